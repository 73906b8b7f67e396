// Context layout shared by the stage sources.
#pragma once
#include "common.cuh"

namespace fv3b {
constexpr int NWS = 40;   // 3-D scratch fields in the workspace
// the last workspace field is the second scratch of the del-n ping-pong
// (delnflux_nosg); no stage uses it for anything else
constexpr int WS_DELN_ALT = NWS - 1;
constexpr int NCOL = 32;  // per-level column arrays
constexpr int MAXLEV = 128;

// indices of the per-level columns in ctx->col
enum ColumnId {
  COL_NORD = 0, COL_NORD_V, COL_NORD_W, COL_NORD_T, COL_DAMP_VT, COL_DAMP_W, COL_DAMP_T, COL_D2_DIVG,
  COL_D_CON, COL_KE_BG, COL_DAMP4_VT_C, COL_DAMP4_W_C, COL_DAMP4_VT, COL_DAMP4_T, COL_DAMP_VT_DZ, COL_SPARE1,
  // acoustic driver columns (AcousticDynamics.__init__): reference layer
  // thickness, cubic-spline constants of UpdateHeightOnDGrid, Rayleigh
  // damping factors
  COL_DP_REF = 16, COL_SPLINE_GK, COL_SPLINE_BETA, COL_SPLINE_GAMMA, COL_RF, COL_RF_DM, COL_DP_RAY
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
  // power-of-two range scales of the del-n passes (1 in double builds) and
  // dd8 divided by area_scale_c^nonzero_nord
  double area_scale = 1.0, area_scale_c = 1.0, dd8_scaled = 0.0;
};

// RayleighDamping per-level factors, recomputed when their inputs change
struct RayState {
  bool ready = false;
  double dt = 0, ptop = 0, rf_cutoff = 0, tau = 0;
  double dp[MAXLEV], pfull[MAXLEV];
  int k_rf = 0, k_nudge = 0;
};

struct AcousticState;  // dyn_core.cu
}  // namespace fv3b

struct fv3b_ctx {
  fv3b::Dims d;
  fv3b_metrics m;
  fv3b::real* ws_base = nullptr;
  fv3b::real* ws[fv3b::NWS];
  fv3b::real* col = nullptr;  // [NCOL][MAXLEV] device columns
  fv3b::DswSetup dsw;
  bool dzd_ready = false;
  int dzd_hord_tm = 0;
  fv3b::RayState ray;
  fv3b::AcousticState* acoustic = nullptr;
  // LagrangianToEulerian: ak and bk in FP64 on the device (2 x MAXLEV),
  // set by fv3b_remap_setup
  double* remap_akbk = nullptr;
  int remap_nlev = 0;
  // the saturation adjustment's tables (es and its differences over water
  // and ice), [4][2624] doubles, filled by fv3b_remap_setup
  double* sat_tables = nullptr;
};

namespace fv3b {
// device pointer of per-level column `id`
inline real* colp(fv3b_ctx* c, int id) { return c->col + (size_t)id * MAXLEV; }
}  // namespace fv3b

// frees the acoustic driver's temporaries (dyn_core.cu)
void fv3b_acoustics_release(fv3b_ctx* ctx);

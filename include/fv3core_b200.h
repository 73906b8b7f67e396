/*
 * fv3core_b200 — C ABI of the B200-native acoustic substep.
 *
 * Every entry point replaces one stencil class (or class method) of the
 * reference, fv3core, whose Python interface is cited beside it.  The
 * reference runs one cube tile per MPI rank; here all six tiles live in one
 * device allocation and every call advances all of them.
 *
 * Memory layout (device pointers, FP64 unless stated):
 *   3-D field   double[6][npz+1][n+2h+1][n+2h+1]   (i fastest)
 *   2-D field   double[6][n+2h+1][n+2h+1]
 *   1-D field   double[npz+1]
 * Index (i, j) in a field is the reference's storage index: the compute
 * domain of a tile is i, j in [h, h+n) (cell centres) or [h, h+n] (edges).
 *
 * All calls are asynchronous on the given CUDA stream (cudaStream_t passed
 * as void*), allocate nothing, and return 0 on success or an FV3B_ERR_*
 * code; fv3b_last_error() describes the last failure of the calling thread.
 */
#ifndef FV3CORE_B200_H
#define FV3CORE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  FV3B_OK = 0,
  FV3B_ERR_ARGUMENT = 1,    /* bad size, null pointer or unsupported option */
  FV3B_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  FV3B_ERR_UNSUPPORTED = 3, /* configuration the reference also rejects */
  FV3B_ERR_TIMEOUT = 4      /* a bounded device wait gave up */
};

typedef struct fv3b_grid_dims {
  int32_t npx;    /* compute cells along a tile edge (n) */
  int32_t n_halo; /* halo width h (3) */
  int32_t npz;    /* number of layers */
  int32_t reserved;
} fv3b_grid_dims;

/*
 * Grid metric terms (device pointers, owned by the caller, read only).
 * 2-D fields are [6][n+2h+1][n+2h+1]; the four edge factors are
 * [6][n+1] (index = position along the tile edge).  Replaces the reference's
 * GridData / DampingCoefficients containers (fv3core/utils/grid.py:475-799)
 * plus the legacy spec.grid fields the hot path reads (fC, f0, agrid, bgrid,
 * edge_*, divg_*).
 */
typedef struct fv3b_metrics {
  const double *dx, *dy, *dxa, *dya, *dxc, *dyc;
  const double *rdx, *rdy, *rdxa, *rdya, *rdxc, *rdyc;
  const double *area, *rarea, *rarea_c;
  const double *sin_sg1, *sin_sg2, *sin_sg3, *sin_sg4;
  const double *cos_sg1, *cos_sg2, *cos_sg3, *cos_sg4;
  const double *cosa, *cosa_u, *cosa_v, *cosa_s, *sina_u, *sina_v;
  const double *rsina, *rsin_u, *rsin_v, *rsin2;
  const double *del6_u, *del6_v, *divg_u, *divg_v;
  const double *fC, *f0;
  const double *agrid1, *agrid2, *bgrid1, *bgrid2;
  const double *edge_w, *edge_e, *edge_s, *edge_n;
  double da_min, da_min_c;
} fv3b_metrics;

/* Opaque context: grid sizes, metric pointers and the device workspace
 * (scratch fields) of the stage kernels.  Created once per grid; stage calls
 * allocate nothing. */
typedef struct fv3b_ctx fv3b_ctx;

/* Allocates the workspace (cudaMalloc) on the current device. */
int fv3b_ctx_create(const fv3b_grid_dims* dims, const fv3b_metrics* metrics, fv3b_ctx** out);
int fv3b_ctx_destroy(fv3b_ctx* ctx);

/*
 * CGridShallowWaterDynamics.__call__ (fv3core/stencils/c_sw.py:534-659)
 * including DGrid2AGrid2CGridVectors (fv3core/stencils/d2a2c_vect.py:543-651)
 * and divergence_corner when nord > 0.
 * In: u, v.  In/out: delp, pt, w (cube-corner halos are filled, as in the
 * reference), uc, vc, ua, va, ut, vt, divgd, omga.  Out: delpc, ptc.
 */
int fv3b_c_sw(fv3b_ctx* ctx, double* delp, double* pt, const double* u, const double* v, double* w,
              double* uc, double* vc, double* ua, double* va, double* ut, double* vt, double* divgd,
              double* omga, double dt2, int nord, double* delpc, double* ptc, void* stream);

/*
 * D-grid shallow-water namelist (DGridShallowWaterLagrangianDynamicsConfig,
 * fv3core/_config.py:137-160).  Flags are 0/1.
 */
typedef struct fv3b_dsw_config {
  double dddmp, d2_bg, d2_bg_k1, d2_bg_k2, d4_bg, ke_bg, d_con, vtdm4, d_ext;
  int32_t nord, n_sponge, grid_type;
  int32_t hord_dp, hord_tm, hord_mt, hord_vt;
  int32_t do_vort_damp, hydrostatic, do_f3d, do_skeb, inline_q, convert_ke;
} fv3b_dsw_config;

/*
 * DGridShallowWaterLagrangianDynamics.__init__ (fv3core/stencils/d_sw.py:611-841):
 * derives the per-level damping columns (get_column_namelist, d_sw.py:512-563)
 * and damping coefficients and stores them in the context.  Rejects the
 * options the reference rejects (grid_type >= 3, inline_q, d_ext > 0,
 * damping columns <= 1e-5) with FV3B_ERR_UNSUPPORTED.
 */
int fv3b_d_sw_setup(fv3b_ctx* ctx, const fv3b_dsw_config* config);

/*
 * DGridShallowWaterLagrangianDynamics.__call__ (fv3core/stencils/d_sw.py:843-1131):
 * FiniteVolumeFluxPrep, five FiniteVolumeTransport calls with del-n damping,
 * kinetic-energy and vorticity terms, DivergenceDamping (with a2b_ord4) and
 * the heat source.  Argument meaning as in the reference; all arrays are
 * 3-D device fields.
 */
int fv3b_d_sw(fv3b_ctx* ctx, double* delpc, double* delp, double* ptc, double* pt, double* u, double* v,
              double* w, double* uc, double* vc, const double* ua, const double* va, double* divgd,
              double* mfx, double* mfy, double* cx, double* cy, double* crx, double* cry, double* xfx,
              double* yfx, double* q_con, const double* zh, double* heat_source, double* diss_est,
              double dt, void* stream);

/* Description of the last error raised on the calling host thread. */
const char* fv3b_last_error(void);

/* Library version string. */
const char* fv3b_version(void);

/*
 * RiemannSolverC.__call__  (fv3core/stencils/riem_solver_c.py:106-165,
 * with Sim1Solver, fv3core/stencils/sim1_solver.py:11-175).
 * Columns i, j in [h-1, h+n] of all tiles, interface levels 0..npz.
 * In: cappa, hs (2-D), ws (2-D), ptc, q_con, delpc, w3.  In/out: gz
 * (heights in, geopotential out).  Out: pef.
 */
int fv3b_riem_solver_c(const fv3b_grid_dims* dims, double dt2, double ptop, double p_fac,
                       const double* cappa, const double* hs, const double* ws,
                       const double* ptc, const double* q_con, const double* delpc,
                       double* gz, double* pef, const double* w3, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FV3CORE_B200_H */

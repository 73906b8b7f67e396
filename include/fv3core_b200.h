/*
 * fv3core_b200 — C ABI of the B200-native acoustic substep.
 *
 * Every entry point replaces one stencil class (or class method) of the
 * reference, fv3core, whose Python interface is cited beside it.  The
 * reference runs one cube tile per MPI rank; here all six tiles live in one
 * device allocation and every call advances all of them.
 *
 * Memory layout (device pointers of fv3b_real, defined below):
 *   3-D field   fv3b_real[6][npz+1][n+2h+1][n+2h+1]   (i fastest)
 *   2-D field   fv3b_real[6][n+2h+1][n+2h+1]
 *   1-D field   fv3b_real[npz+1]
 * Index (i, j) in a field is the reference's storage index: the compute
 * domain of a tile is i, j in [h, h+n) (cell centres) or [h, h+n] (edges).
 *
 * Stage calls are asynchronous on the given CUDA stream (cudaStream_t passed
 * as void*), allocate nothing, and return 0 on success or an FV3B_ERR_*
 * code; fv3b_last_error() describes the last failure of the calling thread.
 * Only fv3b_ctx_create and the *_setup calls allocate or synchronise.
 */
#ifndef FV3CORE_B200_H
#define FV3CORE_B200_H

#include <stdint.h>

/*
 * Field element type.  libfv3core_b200.so is the FP64 build (fv3b_real =
 * double).  libfv3core_b200_f32.so is the mixed-precision build of the same
 * sources (compile with FV3B_REAL_T=float to use it): fields and metric
 * terms are FP32 in memory and the bulk arithmetic is FP32, while the
 * Riemann solvers' column solves, the pe/peln/pk log-pressure integration
 * and the delp column sums run in FP64.  Scalars, configuration structs and
 * host arrays are double in both builds.
 */
#ifndef FV3B_REAL_T
#define FV3B_REAL_T double
#endif
typedef FV3B_REAL_T fv3b_real;

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
 * [6][n+1] (index = position along the tile edge); a2b_extrap is [6][4][3].  Replaces the reference's
 * GridData / DampingCoefficients containers (fv3core/utils/grid.py:475-799)
 * plus the legacy spec.grid fields the hot path reads (fC, f0, agrid, bgrid,
 * edge_*, divg_*).
 */
typedef struct fv3b_metrics {
  const fv3b_real *dx, *dy, *dxa, *dya, *dxc, *dyc;
  const fv3b_real *rdx, *rdy, *rdxa, *rdya, *rdxc, *rdyc;
  const fv3b_real *area, *rarea, *rarea_c;
  const fv3b_real *sin_sg1, *sin_sg2, *sin_sg3, *sin_sg4;
  const fv3b_real *cos_sg1, *cos_sg2, *cos_sg3, *cos_sg4;
  const fv3b_real *cosa, *cosa_u, *cosa_v, *cosa_s, *sina_u, *sina_v;
  const fv3b_real *rsina, *rsin_u, *rsin_v, *rsin2;
  const fv3b_real *del6_u, *del6_v, *divg_u, *divg_v;
  const fv3b_real *fC, *f0;
  const fv3b_real *agrid1, *agrid2, *bgrid1, *bgrid2;
  const fv3b_real *edge_w, *edge_e, *edge_s, *edge_n;
  /* [6][4][3]: x1 / (x2 - x1) of a2b_ord4's cube-corner extrapolations
   * (a2b_ord4.py:38-57), corners (is, js), (ie+1, js), (ie+1, je+1),
   * (is, je+1), three extrapolations each in the reference's order */
  const fv3b_real* a2b_extrap;
  double da_min, da_min_c;
} fv3b_metrics;

/* Opaque context: grid sizes, metric pointers and the device workspace
 * (scratch fields) of the stage kernels.  Created once per grid; stage calls
 * allocate nothing. */
typedef struct fv3b_ctx fv3b_ctx;

/* Allocates the workspace (cudaMalloc) on the current device. */
int fv3b_ctx_create(const fv3b_grid_dims* dims, const fv3b_metrics* metrics, fv3b_ctx** out);

/*
 * A context for an ensemble of `members` cubes of the same grid, advanced
 * together: every array of the context's calls holds 6 x members tile slots
 * (member m owns tiles 6m .. 6m+5, i.e. fields fv3b_real[6 x members][npz+1]
 * [n+2h+1][n+2h+1]), including the metric terms, which the caller repeats
 * for every member.  Each stage call then advances all members in one
 * launch per kernel; halo updates stay within a member.  The reference has
 * no counterpart (it runs one cube per process); it replaces running
 * members one at a time, one context each.  The adjoint entry
 * points serve single cubes only.
 */
int fv3b_ctx_create_batched(const fv3b_grid_dims* dims, const fv3b_metrics* metrics, int members, fv3b_ctx** out);
int fv3b_ctx_destroy(fv3b_ctx* ctx);

/*
 * CGridShallowWaterDynamics.__call__ (fv3core/stencils/c_sw.py:534-659)
 * including DGrid2AGrid2CGridVectors (fv3core/stencils/d2a2c_vect.py:543-651)
 * and divergence_corner when nord > 0.
 * In: u, v.  In/out: delp, pt, w (cube-corner halos are filled, as in the
 * reference), uc, vc, ua, va, ut, vt, divgd, omga.  Out: delpc, ptc.
 */
int fv3b_c_sw(fv3b_ctx* ctx, fv3b_real* delp, fv3b_real* pt, const fv3b_real* u, const fv3b_real* v, fv3b_real* w,
              fv3b_real* uc, fv3b_real* vc, fv3b_real* ua, fv3b_real* va, fv3b_real* ut, fv3b_real* vt, fv3b_real* divgd,
              fv3b_real* omga, double dt2, int nord, fv3b_real* delpc, fv3b_real* ptc, void* stream);

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
int fv3b_d_sw(fv3b_ctx* ctx, fv3b_real* delpc, fv3b_real* delp, fv3b_real* ptc, fv3b_real* pt, fv3b_real* u, fv3b_real* v,
              fv3b_real* w, fv3b_real* uc, fv3b_real* vc, const fv3b_real* ua, const fv3b_real* va, fv3b_real* divgd,
              fv3b_real* mfx, fv3b_real* mfy, fv3b_real* cx, fv3b_real* cy, fv3b_real* crx, fv3b_real* cry, fv3b_real* xfx,
              fv3b_real* yfx, fv3b_real* q_con, const fv3b_real* zh, fv3b_real* heat_source, fv3b_real* diss_est,
              double dt, void* stream);

/* Description of the last error raised on the calling host thread. */
const char* fv3b_last_error(void);

/* Library version string. */
const char* fv3b_version(void);

/* Number of kernel launches this library has issued since it was loaded
 * (diagnostic; all host threads). */
long long fv3b_launch_count(void);

/* Thread-block shapes of the stencil kernels: box kernels get box_x * box_y
 * threads (box_x a multiple of 32, at most 1024 threads), column kernels col
 * threads (a multiple of 32).  Process-wide; results do not depend on it.
 * fv3core_b200.autotune picks it by timing. */
int fv3b_set_launch_shape(int box_x, int box_y, int col);
void fv3b_get_launch_shape(int* box_x, int* box_y, int* col);

/*
 * RiemannSolverC.__call__  (fv3core/stencils/riem_solver_c.py:106-165,
 * with Sim1Solver, fv3core/stencils/sim1_solver.py:11-175).
 * Columns i, j in [h-1, h+n] of all tiles, interface levels 0..npz.
 * In: cappa, hs (2-D), ws (2-D), ptc, q_con, delpc, w3.  In/out: gz
 * (heights in, geopotential out).  Out: pef.
 */
int fv3b_riem_solver_c(const fv3b_grid_dims* dims, double dt2, double ptop, double p_fac,
                       const fv3b_real* cappa, const fv3b_real* hs, const fv3b_real* ws,
                       const fv3b_real* ptc, const fv3b_real* q_con, const fv3b_real* delpc,
                       fv3b_real* gz, fv3b_real* pef, const fv3b_real* w3, void* stream);

/*
 * RiemannSolver3.__call__ (fv3core/stencils/riem_solver3.py:145-242) with
 * a_imp > 0.999, beta = 0, use_logp = False: compute-domain columns,
 * interface levels 0..npz.  In: cappa, zs (2-D), wsd (2-D), q_con, delp, pt.
 * In/out: delz, zh, w, pk3 (levels 0..npz of the compute domain).  Out: ppe
 * (nonhydrostatic pressure perturbation); when last_call != 0 also pe, pk
 * and peln.
 */
int fv3b_riem_solver3(const fv3b_grid_dims* dims, int last_call, double dt, double ptop, double p_fac,
                      const fv3b_real* cappa, const fv3b_real* zs, const fv3b_real* wsd, fv3b_real* delz,
                      const fv3b_real* q_con, const fv3b_real* delp, const fv3b_real* pt, fv3b_real* zh, fv3b_real* pe,
                      fv3b_real* ppe, fv3b_real* pk3, fv3b_real* pk, fv3b_real* peln, fv3b_real* w, void* stream);

/*
 * Adjoint of fv3b_riem_solver3's column solve (no reference counterpart: the
 * reference has no derivatives).  For the compute-domain columns, given the
 * solver's inputs w, zh, delp, pt, wsd (held fixed: cappa, q_con) and the
 * cotangents gw_out of the new w and gdz_out of the new delz (layer levels
 * 0..npz-1), writes the gradients g_w, g_delp, g_pt (layers), g_zh
 * (interfaces 0..npz) and g_wsd (2-D, the surface w) of <gw_out, w_new> +
 * <gdz_out, delz_new>.  The branch of the pressure floor is the forward's.
 * Needs npz >= 3.  It recomputes the forward column in the thread's local
 * memory: correct, not yet fast.
 */
int fv3b_riem_solver3_adjoint(const fv3b_grid_dims* dims, double dt, double ptop, double p_fac,
                              const fv3b_real* cappa, const fv3b_real* wsd, const fv3b_real* q_con,
                              const fv3b_real* delp, const fv3b_real* pt, const fv3b_real* zh, const fv3b_real* w,
                              const fv3b_real* gw_out, const fv3b_real* gdz_out, fv3b_real* g_w, fv3b_real* g_zh,
                              fv3b_real* g_delp, fv3b_real* g_pt, fv3b_real* g_wsd, void* stream);

/*
 * Adjoint of fv3b_riem_solver_c (no reference counterpart).  For the columns
 * is-1..ie+1 x js-1..je+1, given the solver's inputs w3, gz, delpc, ptc, ws
 * (held fixed: cappa, q_con, hs) and the cotangents gpef_out, ggz_out
 * of its outputs pef and gz (interfaces 0..npz), writes the gradients g_w3,
 * g_delpc, g_ptc (layers), g_gz (the input heights, interfaces) and g_ws
 * (2-D, the surface w).  Same conditions as fv3b_riem_solver3_adjoint.
 */
int fv3b_riem_solver_c_adjoint(const fv3b_grid_dims* dims, double dt2, double ptop, double p_fac,
                               const fv3b_real* cappa, const fv3b_real* ws, const fv3b_real* q_con,
                               const fv3b_real* delpc, const fv3b_real* ptc, const fv3b_real* gz, const fv3b_real* w3,
                               const fv3b_real* gpef_out, const fv3b_real* ggz_out, fv3b_real* g_w3,
                               fv3b_real* g_gz, fv3b_real* g_delpc, fv3b_real* g_ptc, fv3b_real* g_ws, void* stream);

/*
 * UpdateGeopotentialHeightOnCGrid.__call__ (fv3core/stencils/updatedzc.py:123-163).
 * dp_ref: device [npz+1] reference layer thickness; zs, ws: 2-D.
 * In: ut, vt.  In/out: gz (interface heights).  Out: ws.
 */
int fv3b_update_dz_c(fv3b_ctx* ctx, const fv3b_real* dp_ref, const fv3b_real* zs, const fv3b_real* ut, const fv3b_real* vt,
                     fv3b_real* gz, fv3b_real* ws, double dt, void* stream);

/*
 * Adjoint of fv3b_update_dz_c (no reference counterpart).  gz is the input
 * heights of the forward call (before it updated them), ut and vt its
 * fluxes; g_gz_out and g_ws are the cotangents of the new gz (3-D) and ws
 * (2-D).  Writes, on every point, the gradients g_gz (of the input heights,
 * the pass-through outside the updated box included), g_ut and g_vt.
 * dp_ref, zs and the areas are held fixed; the upwind choices and the DZ_MIN
 * floor are the forward's.  Uses the context's workspace.
 */
int fv3b_update_dz_c_adjoint(fv3b_ctx* ctx, const fv3b_real* dp_ref, const fv3b_real* ut, const fv3b_real* vt,
                             const fv3b_real* gz, const fv3b_real* g_gz_out, const fv3b_real* g_ws, fv3b_real* g_gz,
                             fv3b_real* g_ut, fv3b_real* g_vt, double dt, void* stream);

/*
 * UpdateHeightOnDGrid.__init__ (fv3core/stencils/updatedzd.py:189-320):
 * dp_ref_host is the host [npz+1] reference layer thickness (dp0), hord_tm
 * the PPM order of the height transport.  Needs
 * fv3b_d_sw_setup first (the damping column namelist).  Synchronous.
 */
int fv3b_update_dz_d_setup(fv3b_ctx* ctx, const double* dp_ref_host, int hord_tm);

/*
 * UpdateHeightOnDGrid.__call__ (fv3core/stencils/updatedzd.py:323-393).
 * In: zs (2-D), crx, cry, xfx, yfx.  In/out: zh.  Out: wsd (2-D).
 */
int fv3b_update_dz_d(fv3b_ctx* ctx, const fv3b_real* zs, fv3b_real* zh, const fv3b_real* crx, const fv3b_real* cry,
                     const fv3b_real* xfx, const fv3b_real* yfx, fv3b_real* wsd, double dt, void* stream);

/* p_grad_c_stencil (fv3core/stencils/dyn_core.py:101-145), nonhydrostatic. */
int fv3b_p_grad_c(fv3b_ctx* ctx, fv3b_real* uc, fv3b_real* vc, const fv3b_real* delpc, const fv3b_real* pkc,
                  const fv3b_real* gz, double dt2, void* stream);

/*
 * Adjoint of fv3b_p_grad_c (no reference counterpart).  Given the inputs
 * delpc, pkc, gz of the forward call and the cotangents gu, gv of the new
 * uc, vc, writes the gradients g_delpc, g_pkc, g_gz of <gu, uc_new> +
 * <gv, vc_new> on [is-1, ie+1] x [js-1, je+1] x levels 0..npz (g_delpc is
 * 0 on level npz); the caller zeroes the points outside that box.  The
 * gradients of uc and vc are gu and gv themselves.
 */
int fv3b_p_grad_c_adjoint(fv3b_ctx* ctx, const fv3b_real* delpc, const fv3b_real* pkc, const fv3b_real* gz,
                          const fv3b_real* gu, const fv3b_real* gv, fv3b_real* g_delpc, fv3b_real* g_pkc,
                          fv3b_real* g_gz, double dt2, void* stream);

/*
 * NonHydrostaticPressureGradient.__call__ (fv3core/stencils/nh_p_grad.py:147-206).
 * pp, pk3 and gz are replaced by their B-grid values, as in the reference.
 */
int fv3b_nh_p_grad(fv3b_ctx* ctx, fv3b_real* u, fv3b_real* v, fv3b_real* pp, fv3b_real* gz, fv3b_real* pk3, fv3b_real* delp,
                   double dt, double ptop, double akap, void* stream);

/*
 * Adjoint of fv3b_nh_p_grad (no reference counterpart).  pp, gz, pk3, delp
 * are the forward call's inputs (before it replaced pp, gz, pk3 by their
 * B-grid values); gu, gv, gpp, ggz, gpk3 the cotangents of its outputs u, v,
 * pp, gz, pk3.  Writes, on every point, the gradients g_u, g_v, g_pp, g_gz,
 * g_pk3 (pass-through outside what the stage writes included) and g_delp.
 * Uses the context's workspace.
 */
int fv3b_nh_p_grad_adjoint(fv3b_ctx* ctx, const fv3b_real* pp, const fv3b_real* gz, const fv3b_real* pk3,
                           const fv3b_real* delp, const fv3b_real* gu, const fv3b_real* gv, const fv3b_real* gpp,
                           const fv3b_real* ggz, const fv3b_real* gpk3, fv3b_real* g_u, fv3b_real* g_v,
                           fv3b_real* g_pp, fv3b_real* g_gz, fv3b_real* g_pk3, fv3b_real* g_delp, double dt,
                           double ptop, double akap, void* stream);

/* edge_pe (fv3core/stencils/pe_halo.py:6-33). */
int fv3b_edge_pe(fv3b_ctx* ctx, fv3b_real* pe, const fv3b_real* delp, double ptop, void* stream);

/* PK3Halo.__call__ (fv3core/stencils/pk3_halo.py:36-68). */
int fv3b_pk3_halo(fv3b_ctx* ctx, fv3b_real* pk3, const fv3b_real* delp, double ptop, double akap, void* stream);

/*
 * Adjoints of fv3b_edge_pe and fv3b_pk3_halo (no reference counterpart).
 * g_pe / g_pk3 hold the cotangent of the new field on entry and that of the
 * old field on return (zero where the stage overwrote it); g_delp is
 * overwritten on every point.  pk3's needs npz <= 127.
 */
int fv3b_edge_pe_adjoint(fv3b_ctx* ctx, fv3b_real* g_pe, fv3b_real* g_delp, void* stream);
int fv3b_pk3_halo_adjoint(fv3b_ctx* ctx, const fv3b_real* delp, fv3b_real* g_pk3, fv3b_real* g_delp, double ptop,
                          double akap, void* stream);

/*
 * RayleighDamping.__call__ (fv3core/stencils/ray_fast.py:169-192); the
 * constructor arguments rf_cutoff, tau, hydrostatic are passed per call.
 * dp and pfull are HOST arrays of npz values (the reference's K fields);
 * factors are re-uploaded (synchronously) only when they change.
 */
int fv3b_ray_fast(fv3b_ctx* ctx, fv3b_real* u, fv3b_real* v, fv3b_real* w, const double* dp, const double* pfull,
                  double dt, double ptop, double rf_cutoff, double tau, int hydrostatic, void* stream);

/*
 * Adjoint of fv3b_ray_fast (no reference counterpart), in place on the
 * cotangents gu, gv, gw of the new winds.  Uses the damping constants of
 * the last fv3b_ray_fast call on this context, whose arguments these must
 * match (FV3B_ERR_ARGUMENT otherwise).
 */
int fv3b_ray_fast_adjoint(fv3b_ctx* ctx, fv3b_real* gu, fv3b_real* gv, fv3b_real* gw, const double* dp,
                          const double* pfull, double dt, double ptop, double rf_cutoff, double tau, int hydrostatic,
                          void* stream);

/* HyperdiffusionDamping.__call__ (fv3core/stencils/del2cubed.py:152-181). */
int fv3b_del2cubed(fv3b_ctx* ctx, fv3b_real* qdel, double cd, int nmax, void* stream);

/*
 * Adjoint of fv3b_del2cubed (no reference counterpart), in place: gq holds
 * the cotangent of the filtered field on entry and that of the field before
 * the filter on return.  Uses the context's workspace.
 */
int fv3b_del2cubed_adjoint(fv3b_ctx* ctx, fv3b_real* gq, double cd, int nmax, void* stream);

/* compute_pkz_tempadjust (fv3core/stencils/temperature_adjust.py:8-44) on
 * levels [0, nk_heat). */
int fv3b_pkz_tempadjust(fv3b_ctx* ctx, const fv3b_real* delp, const fv3b_real* delz, const fv3b_real* cappa,
                        const fv3b_real* heat_source, fv3b_real* pt, fv3b_real* pkz, double delt_time_factor, int nk_heat,
                        void* stream);

/*
 * Adjoint of fv3b_pkz_tempadjust (no reference counterpart).  delp, delz,
 * cappa, heat_source, pt: the forward call's inputs.  g_pt, g_pkz: the
 * cotangents of the new pt, pkz on entry, of the old ones on return.
 * g_delp, g_delz, g_heat: overwritten on every point.  cappa is held fixed.
 */
int fv3b_pkz_tempadjust_adjoint(fv3b_ctx* ctx, const fv3b_real* delp, const fv3b_real* delz, const fv3b_real* cappa,
                                const fv3b_real* heat_source, const fv3b_real* pt, fv3b_real* g_pt, fv3b_real* g_pkz,
                                fv3b_real* g_delp, fv3b_real* g_delz, fv3b_real* g_heat, double delt_time_factor,
                                int nk_heat, void* stream);

/*
 * Halo updates, replacing fv3gfs-util's HaloUpdater.update /
 * CubedSphereCommunicator.synchronize_vector_interfaces as the reference's
 * AcousticDynamics._HaloUpdaters use them (fv3core/stencils/dyn_core.py:216-286).
 * All six tiles are in one allocation, so an update is an on-device gather.
 * stagger: 1 = cell centres, 0 = cell corners.  grid: 0 = D-grid (u, v),
 * 1 = C-grid (uc, vc).  nlev: levels to update (npz for Z_DIM fields,
 * npz+1 for Z_INTERFACE_DIM fields).
 */
int fv3b_halo_update_scalar(fv3b_ctx* ctx, fv3b_real* field, int stagger, int n_halo, int nlev, void* stream);
int fv3b_halo_update_vector(fv3b_ctx* ctx, fv3b_real* x, fv3b_real* y, int grid, int nlev, void* stream);
int fv3b_synchronize_vector_interfaces(fv3b_ctx* ctx, fv3b_real* u, fv3b_real* v, int nlev, void* stream);

/*
 * Adjoints of the three halo calls above (no reference counterpart), in
 * place: on entry the arrays hold the cotangents of the updated fields, on
 * return those of the fields before the update (each halo point's
 * cotangent added into its source, rotated like the forward copy, and the
 * halo point zeroed).  Same arguments and conditions as the forward calls.
 */
int fv3b_halo_update_scalar_adjoint(fv3b_ctx* ctx, fv3b_real* g, int stagger, int n_halo, int nlev, void* stream);
int fv3b_halo_update_vector_adjoint(fv3b_ctx* ctx, fv3b_real* gx, fv3b_real* gy, int grid, int nlev, void* stream);
int fv3b_synchronize_vector_interfaces_adjoint(fv3b_ctx* ctx, fv3b_real* gu, fv3b_real* gv, int nlev,
                                               void* stream);

/*
 * AcousticDynamicsConfig (fv3core/_config.py:164-212) without the nested
 * RiemannConfig / D-grid config (p_fac comes from the Riemann config; the
 * D-grid namelist is passed separately).  Flags are 0/1.
 */
typedef struct fv3b_acoustic_config {
  double tau, delt_max, rf_cutoff, p_fac;
  int32_t k_split, n_split, rf_fast, breed_vortex_inline, use_old_omega, reserved;
} fv3b_acoustic_config;

/*
 * The dycore state fields AcousticDynamics.__call__ reads and writes
 * (fv3core/stencils/dyn_core.py:479-761), as device pointers in the layout
 * above; phis and wsd are 2-D.  mdt, n_map, akap, ptop, ks are the state's
 * scalars.
 */
typedef struct fv3b_dycore_state {
  fv3b_real *u, *v, *w, *delz, *delp, *pt, *pe, *pk, *phis, *wsd, *omga, *ua, *va, *uc, *vc;
  fv3b_real *mfxd, *mfyd, *cxd, *cyd, *pkz, *peln, *q_con, *diss_estd, *cappa;
  double mdt, akap, ptop;
  int32_t n_map, ks;
} fv3b_dycore_state;

/*
 * AcousticDynamics.__init__ (fv3core/stencils/dyn_core.py:288-477): D-grid
 * setup, reference layer thickness dp_ref from ak/bk, zs = phis/g, spline
 * constants, and the substep temporaries (gz, zh, pkc, pk3, ut, vt, divgd,
 * heat_source, crx, cry, xfx, yfx, delpc, ptc, ws3), which persist between
 * calls as the reference's instance storages do.  ak, bk, pfull: HOST
 * arrays of npz+1, npz+1, npz values; phis: device 2-D field.  Allocates
 * (cudaMalloc) and synchronises.  Rejects what the reference rejects
 * (d_ext != 0, beta != 0, use_logp, hydrostatic).
 */
int fv3b_acoustics_setup(fv3b_ctx* ctx, const fv3b_acoustic_config* config, const fv3b_dsw_config* dsw,
                         const double* ak, const double* bk, const double* pfull, const fv3b_real* phis);

/*
 * AcousticDynamics.__call__ (fv3core/stencils/dyn_core.py:479-761): the
 * n_split acoustic substeps (c_sw, updatedzc, riem_solver_c, p_grad_c,
 * d_sw, updatedzd, riem_solver3, pe/pk3 halos, nh_p_grad, ray_fast, halo
 * updates) and the closing del2cubed / temperature adjustment.
 */
int fv3b_acoustics(fv3b_ctx* ctx, const fv3b_dycore_state* state, void* stream);

/*
 * FiniteVolumeTransport as an object (fv3core/stencils/fvtp2d.py:151-247,
 * constructor FiniteVolumeTransport(stencil_factory, grid_data,
 * damping_coefficients, grid_type, hord, nord=None, damp_c=None)).  hord is
 * the PPM order (5, 6, 7, or 8 for the ord-8 limiter of tracer transport);
 * nord and damp_c are HOST per-level columns of n >= npz values (both NULL
 * for no del-n damping), turned into the DelnFlux coefficients
 * (damp_c * da_min)^(nord + 1) (delnflux.py:24-26, 907-962).  Allocates the
 * device columns (cudaMalloc) and synchronises.  Rejects damp_c columns
 * that are small only on some levels (FV3B_ERR_UNSUPPORTED), as DelnFlux
 * does.  Lives until fv3b_transport_destroy; belongs to ctx.
 */
typedef struct fv3b_transport fv3b_transport;
int fv3b_transport_create(fv3b_ctx* ctx, int hord, const double* nord, const double* damp_c, int n,
                          fv3b_transport** out);
int fv3b_transport_destroy(fv3b_transport* transport);

/*
 * FiniteVolumeTransport.__call__ (fv3core/stencils/fvtp2d.py:249-362):
 * q_x_flux, q_y_flux = the Lin-Rood fluxes of q from the Courant numbers
 * crx, cry and the area fluxes; x/y_mass_flux (NULL: the area fluxes) weight
 * the final fluxes; mass (NULL allowed without damping) weights the del-n
 * damping.  q's 3x3 cube-corner halo blocks are overwritten with their
 * x-direction copies, as the reference's CopiedCorners base is
 * (corners.py:64-117); its y-direction copies are read on the fly.
 */
int fv3b_fvtp2d(const fv3b_transport* transport, fv3b_real* q, const fv3b_real* crx, const fv3b_real* cry,
                const fv3b_real* x_area_flux, const fv3b_real* y_area_flux, fv3b_real* q_x_flux,
                fv3b_real* q_y_flux, const fv3b_real* x_mass_flux, const fv3b_real* y_mass_flux,
                const fv3b_real* mass, void* stream);

/*
 * XPiecewiseParabolic.__call__ (axis 0; fv3core/stencils/xppm.py:283-347)
 * and YPiecewiseParabolic.__call__ (axis 1; yppm.py): flux = the mean of q
 * advected through each interface for Courant number c, order iord (5, 6, 7
 * or 8), over the box [i0, i0+ni) x [j0, j0+nj) x [k0, k0+nk) (the
 * reference's origin and domain).  The tile-edge rules apply at the tile's
 * compute-domain edges, as the reference's i_start / i_end externals place
 * them.  The box plus three points before and two after along the axis
 * must lie inside the storage.  dxa / dya are the context's.
 */
int fv3b_ppm_flux(fv3b_ctx* ctx, int axis, int iord, const fv3b_real* q, const fv3b_real* c, fv3b_real* flux,
                  int i0, int j0, int k0, int ni, int nj, int nk, void* stream);

/*
 * TracerAdvection.__call__ (fv3core/stencils/tracer_2d_1l.py:199-300),
 * constructed with the given transport (hord_tr, no damping; fv_dynamics.py
 * 301-309): area fluxes from the accumulated Courant numbers cxd, cyd; the
 * fixed three sub-steps (cmax = 2), cxd, cyd, mfxd, mfyd scaled by 1/3 in
 * place; each sub-step adjusts the pressure thickness by the mass-flux
 * divergence and transports and re-weights every tracer, with tracer halo
 * updates in between.  tracers: HOST array of ntracers device pointers
 * (3-D fields), updated in place.  dp1 serves as one of the two pressure
 * thickness buffers and holds the second sub-step's value afterwards, as
 * the reference's does.  mdt is unused, as in the reference.
 */
int fv3b_tracer_advection(const fv3b_transport* transport, int ntracers, fv3b_real* const* tracers,
                          fv3b_real* dp1, fv3b_real* mfxd, fv3b_real* mfyd, fv3b_real* cxd, fv3b_real* cyd,
                          double mdt, void* stream);

/*
 * compute_preamble of DynamicalCore.step_dynamics (fv3core/stencils/
 * fv_dynamics.py:54-106): fv_setup with moist_phys and nwat = 6
 * (moist_cv.py:197-228: cvm, q_con, dp1 = zvir * qvapor, cappa, pkz) followed
 * by pt_adjust (fv_dynamics.py:32-34), in one pass over the compute domain
 * and the npz layers.  Water species, delp, delz in; q_con, cvm, pkz,
 * cappa, dp1 out; pt in and out.
 */
int fv3b_compute_preamble(fv3b_ctx* ctx, const fv3b_real* qvapor, const fv3b_real* qliquid, const fv3b_real* qrain,
                          const fv3b_real* qsnow, const fv3b_real* qice, const fv3b_real* qgraupel,
                          fv3b_real* q_con, fv3b_real* cvm, fv3b_real* pkz, fv3b_real* pt, fv3b_real* cappa,
                          const fv3b_real* delp, const fv3b_real* delz, fv3b_real* dp1, void* stream);

/*
 * post_remap of DynamicalCore.step_dynamics (fv_dynamics.py:109-133) for the
 * nonhydrostatic dynamics: set_omega (omga = delp / delz * w, fv_dynamics.py
 * 37-39) and, when nf_omega > 0, the halo update of omga and nf_omega del-2
 * passes (HyperdiffusionDamping) with coefficient 0.18 da_min.
 */
int fv3b_post_remap(fv3b_ctx* ctx, const fv3b_real* delp, const fv3b_real* delz, const fv3b_real* w,
                    fv3b_real* omga, int nf_omega, void* stream);

/*
 * AdjustNegativeTracerMixingRatio.__call__ (fv3core/stencils/neg_adj3.py
 * 293-372), the first half of wrapup (fv_dynamics.py:136-169): fix_neg_water,
 * fillq on graupel and rain, fix_water_vapor_down and fix_neg_cloud on the
 * compute-domain columns.  hydrostatic != 0 is rejected
 * (FV3B_ERR_UNSUPPORTED), as the reference does.  peln is not read (the
 * reference passes it and does not read it either).
 */
int fv3b_adjust_negative_tracers(fv3b_ctx* ctx, fv3b_real* qvapor, fv3b_real* qliquid, fv3b_real* qrain,
                                 fv3b_real* qsnow, fv3b_real* qice, fv3b_real* qgraupel, fv3b_real* qcld,
                                 fv3b_real* pt, const fv3b_real* delp, const fv3b_real* delz,
                                 const fv3b_real* peln, int hydrostatic, void* stream);

/*
 * CubedToLatLon.__call__ (fv3core/stencils/c2l_ord.py:75-141), the second
 * half of wrapup: D-grid winds u, v to A-grid winds ua, va in longitude /
 * latitude components.  order 4: vector halo update of u, v, then
 * ord4_transform on the compute domain; order 2: c2l_ord2 on the compute
 * domain plus one halo row.  a11 .. a22: 2-D device fields of the
 * transformation (the legacy grid's a11 .. a22, fv3core/grid/geometry.py
 * 596-601).
 */
int fv3b_cubed_to_latlon(fv3b_ctx* ctx, fv3b_real* u, fv3b_real* v, const fv3b_real* a11, const fv3b_real* a12,
                         const fv3b_real* a21, const fv3b_real* a22, fv3b_real* ua, fv3b_real* va, int order,
                         void* stream);

/*
 * LagrangianToEulerian.__init__ (fv3core/stencils/remapping.py:210-414):
 * keeps the hybrid coordinate ak, bk (HOST arrays of npz+1 values) on the
 * device in FP64, and on the first call fills the saturation adjustment's
 * tables (saturation vapour pressure over water and ice and their
 * differences at every table index, 84 KB).  Allocates (cudaMalloc) on the
 * first call for a context and synchronises.
 */
int fv3b_remap_setup(fv3b_ctx* ctx, const double* ak, const double* bk);

/*
 * RemappingConfig (fv3core/_config.py:114-125) without the saturation
 * adjustment: the PPM remapping orders (|kord| <= 10; kord_tm < 0, as the
 * reference requires) and fill (0/1, negative-tracer filling after the
 * tracer remap).
 */
typedef struct fv3b_remap_config {
  int32_t kord_tm, kord_tr, kord_wz, kord_mt, fill, reserved;
} fv3b_remap_config;

/*
 * The fields LagrangianToEulerian.__call__ reads and writes, as device
 * pointers: the eight remapped tracers in the reference's order (qvapor,
 * qliquid, qrain, qice, qsnow, qgraupel, qo3mr, qsgs_tke;
 * fv3core/utils/gt4py_utils.py:26-36), the 3-D state fields, ps (2-D,
 * written) and wsd (2-D, the bottom boundary value of w).
 */
typedef struct fv3b_remap_fields {
  fv3b_real* tracers[8];
  fv3b_real *pt, *delp, *delz, *peln, *u, *v, *w, *ua, *va, *cappa, *q_con, *pkz, *pk, *pe, *ps;
  const fv3b_real* wsd;
  /* read only by the saturation adjustment: the cloud fraction (written),
   * dp1 (the reference passes it as the total-energy field) and the surface
   * geopotential hs (2-D) */
  fv3b_real *qcld, *dp1;
  const fv3b_real* hs;
} fv3b_remap_fields;

/*
 * SatAdjustConfig (fv3core/_config.py:85-110): the fast saturation
 * adjustment's namelist.  Flags are 0/1; hydrostatic must be 0.
 */
typedef struct fv3b_sat_adjust_config {
  double sat_adj0, ql_gen, qs_mlt, ql0_max, t_sub, qi_gen, qi_lim, qi0_max, dw_ocean, dw_land, cld_min;
  double tau_i2s, tau_v2l, tau_r2g, tau_l2r, tau_l2v, tau_imlt, tau_smlt;
  int32_t icloud_f, rad_snow, rad_rain, rad_graupel, tintqs, hydrostatic;
} fv3b_sat_adjust_config;

/*
 * LagrangianToEulerian.__call__ (fv3core/stencils/remapping.py:416-628):
 * moist pt and the delz adjustment, the Eulerian pressures ak + bk ps, the
 * PPM remapping (remap_profile.py cs_profile, map_single.py) of pt in log
 * pressure, of the tracers (then fillz) and of w, delz, u and v, moist pkz,
 * the fast saturation adjustment when ``sat`` is not NULL (do_sat_adj;
 * SatAdjust3d, saturation_adjustment.py:544-1024, on levels [kmp, npz),
 * remapping time step mdt, without the total-energy fixer: consv_te 0),
 * and the last-step pt conversion (last_step 1) or the division by pkz
 * (last_step 0).  The remaps run one thread per column, the adjustment one
 * thread per point; both compute in FP64 in both builds.  Requires
 * fv3b_remap_setup.
 */
int fv3b_lagrangian_to_eulerian(fv3b_ctx* ctx, const fv3b_remap_fields* fields, const fv3b_remap_config* config,
                                const fv3b_sat_adjust_config* sat, double ptop, double akap, double zvir,
                                double mdt, int kmp, int last_step, void* stream);

/* Device pointer of one of the substep temporaries by its reference name
 * ("gz", "zh", "pkc", "pk3", "ut", "vt", "divgd", "heat_source", "crx",
 * "cry", "xfx", "yfx", "delpc", "ptc", "ws3", "zs", "dp_ref"), or NULL. */
fv3b_real* fv3b_acoustics_temporary(fv3b_ctx* ctx, const char* name);

/*
 * fv3b_generate_grid: the metric terms of one cube generated on the device,
 * in place of MetricTerms (fv3core/grid/generation.py:66-2137, with
 * gnomonic.py and geometry.py), which the reference computes on the host,
 * one MPI rank per sub-tile, with halo updates between its steps.  Each
 * output value is a closed-form function of the equiangular gnomonic cube
 * (no halo update, no intermediate array, nothing allocated); the values
 * are those of the package's host generator (fv3core_b200/grid.py) to
 * rounding.  Outputs, all FP64 device arrays the caller allocates:
 *   field[f]: FV3B_GRID_NFIELDS 2-D fields, each [6][m][m] with i fastest,
 *     m = n + 2*halo + 1, in this order: dx dy dxa dya dxc dyc rdx rdy rdxa
 *     rdya rdxc rdyc area rarea area_c rarea_c sin_sg1..5 cos_sg1..5 cosa
 *     sina rsina cosa_u cosa_v cosa_s sina_u sina_v rsin_u rsin_v rsin2
 *     del6_u del6_v divg_u divg_v fC f0 agrid1 agrid2 bgrid1 bgrid2 a11 a12
 *     a21 a22;
 *   edge[e]: the A->B edge weights edge_w, edge_e, edge_s, edge_n, [6][n+1];
 *   a2b_extrap: a2b_ord4's cube-corner extrapolation ratios, [6][4][3];
 *   scalars: da_min, da_max (cell areas over the compute domain), da_min_c,
 *     da_max_c (dual cells over the compute corners), [4].
 * lattice: 0 for the equiangular lattice (the package's default grid), 1
 * for the reference's gnomonic_ed (grid_type 0: edge points equally spaced
 * along the edges, fv3core/grid/global_setup.py:42-85).  radius in m,
 * omega in 1/s (Coriolis fC, f0).  Needs 1 <= halo <= 8 and
 * 2*halo <= n <= 4096.  Kernels run on `stream`; the call returns before
 * they finish.
 */
#define FV3B_GRID_NFIELDS 51
typedef struct {
  double* field[FV3B_GRID_NFIELDS];
  double* edge[4];
  double* a2b_extrap;
  double* scalars;
} fv3b_grid_fields;
int fv3b_generate_grid(int n, int halo, int lattice, double radius, double omega, const fv3b_grid_fields* out,
                       void* stream);

/*
 * fv3b_del2cubed_noalloc: no reference counterpart.  The same filter as
 * fv3b_del2cubed (HyperdiffusionDamping, fv3core/stencils/del2cubed.py:152-181)
 * for callers that cannot let the library allocate device memory: it takes
 * no context (fv3b_ctx_create allocates the full stage workspace) and
 * allocates nothing; its scratch is a fixed file-scope device array of
 * 3 x 1,500,000 elements of fv3b_real (36 MB in the FP64 build, 18 MB in the
 * mixed-precision build), reserved on every device that loads the library.
 * Grids with 6*(npz+1)*(npx+2*n_halo+1)^2 above 1,500,000 (larger than
 * C48 L79) are rejected with FV3B_ERR_ARGUMENT.  A call on a stream that is
 * not capturing looks up the scratch's device address (so the address stays
 * valid after a cudaDeviceReset); a call during stream capture uses the
 * address kept by the last uncaptured call on that device, so the first call
 * on a device must come before any stream capture.  The scratch is shared by
 * every caller on a device and keeps the last call's contents (nothing in it
 * needs to start at zero): calls must not overlap in time (issue them on one
 * stream, or order them).  metrics: as for fv3b_ctx_create (del6_u, del6_v
 * and rarea are read).
 */
int fv3b_del2cubed_noalloc(const fv3b_grid_dims* dims, const fv3b_metrics* metrics, fv3b_real* qdel, double cd, int nmax,
                           void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FV3CORE_B200_H */

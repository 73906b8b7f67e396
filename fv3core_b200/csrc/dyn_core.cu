// AcousticDynamics (fv3core/stencils/dyn_core.py:210-761): the acoustic
// substep loop over all six tiles, calling the stage entry points in the
// reference's order.  The halo exchanges that fv3gfs-util runs as MPI
// messages are on-device gathers (halo.cu).  Everything is enqueued on one
// stream; the host never waits inside a call.
#include <math.h>
#include <string.h>

#include <new>
#include <vector>

#include "ctx.cuh"
#include "halo_ops.cuh"
#include "stencil.cuh"

namespace fv3b {

// fill value of the gz and pk3 temporaries (dyn_core.py:333-336); FP32
// holds 1e30 instead of 1e40
constexpr double HUGE_R = sizeof(real) == sizeof(double) ? 1.0e40 : 1.0e30;
constexpr real GRAV_ = RC(9.80665);
constexpr double KAPPA_ = 287.05 / 1004.6;

enum TmpId {
  T_GZ, T_ZH, T_PKC, T_PK3, T_UT, T_VT, T_DIVGD, T_HEAT, T_CRX, T_CRY, T_XFX, T_YFX, T_DELPC, T_PTC, N_TMP3
};
static const char* const TMP_NAMES[N_TMP3] = {"gz",  "zh",  "pkc", "pk3", "ut",  "vt",    "divgd",
                                              "heat_source", "crx", "cry", "xfx", "yfx", "delpc", "ptc"};

struct AcousticState {
  fv3b_acoustic_config cfg;
  real* base = nullptr;
  real* tmp[N_TMP3];
  real *ws3 = nullptr, *zs = nullptr;
  std::vector<double> dp_ref, pfull;
  int nk_heat = 0;
  bool do_del2cubed = false;
  double cd = 0.0;
};

namespace {
__global__ void fill_kernel(real* p, long long n, real v) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

cudaError_t fill(real* p, long long n, real v, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  fill_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, n, v);
  note_launch();
  return cudaGetLastError();
}

// get_nk_heat_dissipation (dyn_core.py:148-163)
int nk_heat_dissipation(const fv3b_dsw_config& c, int npz) {
  if (c.convert_ke || c.vtdm4 > 1.0e-4) return npz;
  if (c.d2_bg_k1 < 1.0e-3) return 0;
  if (c.d2_bg_k2 < 1.0e-3) return 1;
  return 2;
}
}  // namespace
}  // namespace fv3b

using namespace fv3b;

extern "C" int fv3b_acoustics_setup(fv3b_ctx* ctx, const fv3b_acoustic_config* config, const fv3b_dsw_config* dsw,
                                    const double* ak, const double* bk, const double* pfull, const real* phis) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && config && dsw && ak && bk && pfull && phis, "fv3b_acoustics_setup: null argument");
  FV3B_REQUIRE(dsw->d_ext == 0.0, "fv3b_acoustics_setup: d_ext != 0 is not implemented");
  FV3B_REQUIRE(!dsw->hydrostatic, "fv3b_acoustics_setup: only the nonhydrostatic dynamics are implemented");
  FV3B_REQUIRE(config->n_split >= 1 && config->k_split >= 1, "fv3b_acoustics_setup: n_split, k_split >= 1");
  FV3B_REQUIRE(dsw->grid_type < 4, "fv3b_acoustics_setup: grid_type >= 4 is not implemented");
  const Dims d = ctx->d;
  const int nz = d.nz, nk = d.nk;
  int rc = fv3b_d_sw_setup(ctx, dsw);
  if (rc != FV3B_OK) return rc;
  AcousticState* a = ctx->acoustic;
  if (a == nullptr) {
    a = new (std::nothrow) AcousticState();
    FV3B_REQUIRE(a != nullptr, "fv3b_acoustics_setup: out of host memory");
    const size_t n3 = (size_t)d.st * d.nt, n2 = (size_t)d.st2 * d.nt;
    cudaError_t e = cudaMalloc((void**)&a->base, sizeof(real) * (n3 * N_TMP3 + 2 * n2));
    if (e != cudaSuccess) {
      delete a;
      set_last_error("fv3b_acoustics_setup", e);
      return FV3B_ERR_CUDA;
    }
    for (int q = 0; q < N_TMP3; ++q) a->tmp[q] = a->base + n3 * q;
    a->ws3 = a->base + n3 * N_TMP3;
    a->zs = a->ws3 + n2;
    ctx->acoustic = a;
  }
  a->cfg = *config;
  // dp_ref_compute (dyn_core.py:66-77), K part: layer thickness of the
  // reference column; the bottom interface keeps 0
  a->dp_ref.assign(nk, 0.0);
  for (int k = 0; k < nz; ++k) a->dp_ref[k] = ak[k + 1] - ak[k] + (bk[k + 1] - bk[k]) * 1.0e5;
  a->pfull.assign(pfull, pfull + nz);
  rc = fv3b_update_dz_d_setup(ctx, a->dp_ref.data(), dsw->hord_tm);
  if (rc != FV3B_OK) return rc;
  a->nk_heat = nk_heat_dissipation(*dsw, nz);
  a->do_del2cubed = a->nk_heat != 0 && dsw->d_con > 1.0e-5;
  a->cd = 0.2 * ctx->m.da_min;
  // temporaries: zero, gz and pk3 at HUGE_R (dyn_core.py:333-336)
  const size_t n3 = (size_t)d.st * d.nt, n2 = (size_t)d.st2 * d.nt;
  FV3B_CHECK(cudaMemset(a->base, 0, sizeof(real) * (n3 * N_TMP3 + 2 * n2)));
  FV3B_CHECK(fill(a->tmp[T_GZ], (long long)n3, HUGE_R, 0));
  FV3B_CHECK(fill(a->tmp[T_PK3], (long long)n3, HUGE_R, 0));
  // zs = phis * (1 / g) (dp_ref_compute, dyn_core.py:79)
  real* zs = a->zs;
  FV3B_CHECK(launch_columns(0, d.ni, 0, d.nj, 0, [=] __device__(int t, int i, int j) {
    zs[idx2(d, t, i, j)] = phis[idx2(d, t, i, j)] * (RC(1.0) / GRAV_);
  }));
  FV3B_CHECK(cudaDeviceSynchronize());
  return FV3B_OK;
}

extern "C" real* fv3b_acoustics_temporary(fv3b_ctx* ctx, const char* name) {
  if (!ctx || !ctx->acoustic || !name) return nullptr;
  AcousticState* a = ctx->acoustic;
  for (int q = 0; q < N_TMP3; ++q)
    if (strcmp(name, TMP_NAMES[q]) == 0) return a->tmp[q];
  if (strcmp(name, "ws3") == 0) return a->ws3;
  if (strcmp(name, "zs") == 0) return a->zs;
  if (strcmp(name, "dp_ref") == 0) return colp(ctx, COL_DP_REF);
  return nullptr;
}

void fv3b_acoustics_release(fv3b_ctx* ctx) {
  if (ctx && ctx->acoustic) {
    cudaFree(ctx->acoustic->base);
    delete ctx->acoustic;
    ctx->acoustic = nullptr;
  }
}

#define FV3B_CALL(expr)             \
  do {                              \
    int _rc = (expr);               \
    if (_rc != FV3B_OK) return _rc; \
  } while (0)

extern "C" int fv3b_acoustics(fv3b_ctx* ctx, const fv3b_dycore_state* S, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && S, "fv3b_acoustics: null argument");
  FV3B_REQUIRE(ctx->acoustic, "fv3b_acoustics: call fv3b_acoustics_setup first");
  AcousticState* a = ctx->acoustic;
  const fv3b_acoustic_config& cfg = a->cfg;
  const fv3b_dsw_config& dcfg = ctx->dsw.cfg;
  const Dims d = ctx->d;
  const int nz = d.nz, nk = d.nk;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  const int full = d.ni - 1;
  cudaStream_t st = (cudaStream_t)stream;
  fv3b_grid_dims gd{d.n, d.h, d.nz, 0};
  real** T = a->tmp;
  real *gz = T[T_GZ], *zh = T[T_ZH], *pkc = T[T_PKC], *pk3 = T[T_PK3], *ut = T[T_UT], *vt = T[T_VT];
  real *divgd = T[T_DIVGD], *heat = T[T_HEAT], *crx = T[T_CRX], *cry = T[T_CRY], *xfx = T[T_XFX],
         *yfx = T[T_YFX], *delpc = T[T_DELPC], *ptc = T[T_PTC];
  real *ws3 = a->ws3, *zs = a->zs;
  const real* dp_ref = colp(ctx, COL_DP_REF);
  const int n_split = cfg.n_split;
  const double akap = KAPPA_;
  const double dt = S->mdt / n_split;
  const double dt2 = 0.5 * dt;
  const double ptop = S->ptop;

  {
    real* qc[2] = {S->q_con, S->cappa};
    FV3B_CHECK(halo_scalars(d, qc, 2, 1, d.h, nz, st));
    real* dpt[2] = {S->delp, S->pt};
    FV3B_CHECK(halo_scalars(d, dpt, 2, 1, d.h, nz, st));
    FV3B_CHECK(halo_vector(d, S->u, S->v, false, nz, st));
  }
  // zero_data (dyn_core.py:47-63)
  {
    real *mfxd = S->mfxd, *mfyd = S->mfyd, *cxd = S->cxd, *cyd = S->cyd, *diss = S->diss_estd;
    const bool first = S->n_map == 1;
    FV3B_CHECK(launch_box(Box{0, full, 0, full, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      W3(mfxd, i, j) = RC(0.0);
      W3(mfyd, i, j) = RC(0.0);
      W3(cxd, i, j) = RC(0.0);
      W3(cyd, i, j) = RC(0.0);
      if (first && i >= s && i <= e && j >= js && j <= je) W3(diss, i, j) = RC(0.0);
    }));
  }
  for (int it = 0; it < n_split; ++it) {
    const bool remap_step = cfg.breed_vortex_inline || it == n_split - 1;
    FV3B_CHECK(halo_scalars(d, &S->w, 1, 1, d.h, nz, st));
    if (it == 0) {
      // set_gz (dyn_core.py:80-85) on the compute domain
      const real* delz = S->delz;
      FV3B_CHECK(launch_columns(s, e + 1, js, je + 1, st, [=] __device__(int t, int i, int j) {
        idx_t o = idx3(d, t, i, j, nz);
        double g = zs[idx2(d, t, i, j)];  // column sum in double in every build
        gz[o] = static_cast<real>(g);
        for (int k = nz - 1; k >= 0; --k) {
          o -= d.sk;
          g = g - delz[o];
          gz[o] = static_cast<real>(g);
        }
      }));
      FV3B_CHECK(halo_scalars(d, &gz, 1, 1, d.h, nk, st));
    }
    FV3B_CALL(fv3b_c_sw(ctx, S->delp, S->pt, S->u, S->v, S->w, S->uc, S->vc, S->ua, S->va, ut, vt, divgd, S->omga,
                        dt2, dcfg.nord, delpc, ptc, st));
    if (dcfg.nord > 0) FV3B_CHECK(halo_scalars(d, &divgd, 1, 0, d.h, nz, st));
    // copy_stencil on the full domain, every interface
    {
      const real* src = it == 0 ? gz : zh;
      real* dst = it == 0 ? zh : gz;
      FV3B_CHECK(launch_box(Box{0, full, 0, full, 0, nk}, st, [=] __device__(int t, int i, int j, int k) {
        PT_SETUP(d, t, k);
        W3(dst, i, j) = F3(src, i, j);
      }));
    }
    FV3B_CALL(fv3b_update_dz_c(ctx, dp_ref, zs, ut, vt, gz, ws3, dt2, st));
    FV3B_CALL(fv3b_riem_solver_c(&gd, dt2, ptop, cfg.p_fac, S->cappa, S->phis, ws3, ptc, S->q_con, delpc, gz, pkc,
                                 S->omga, st));
    FV3B_CALL(fv3b_p_grad_c(ctx, S->uc, S->vc, delpc, pkc, gz, dt2, st));
    FV3B_CHECK(halo_vector(d, S->uc, S->vc, true, nz, st));
    FV3B_CALL(fv3b_d_sw(ctx, vt, S->delp, ptc, S->pt, S->u, S->v, S->w, S->uc, S->vc, S->ua, S->va, divgd, S->mfxd,
                        S->mfyd, S->cxd, S->cyd, crx, cry, xfx, yfx, S->q_con, zh, heat, S->diss_estd, dt, st));
    {
      real* f3[3] = {S->delp, S->pt, S->q_con};
      FV3B_CHECK(halo_scalars(d, f3, 3, 1, d.h, nz, st));
    }
    FV3B_CALL(fv3b_update_dz_d(ctx, zs, zh, crx, cry, xfx, yfx, S->wsd, dt, st));
    FV3B_CALL(fv3b_riem_solver3(&gd, remap_step ? 1 : 0, dt, ptop, cfg.p_fac, S->cappa, zs, S->wsd, S->delz,
                                S->q_con, S->delp, S->pt, zh, S->pe, pkc, pk3, S->pk, S->peln, S->w, st));
    FV3B_CHECK(halo_scalars(d, &zh, 1, 1, d.h, nk, st));
    FV3B_CHECK(halo_scalars(d, &pkc, 1, 1, 2, nk, st));
    if (remap_step) FV3B_CALL(fv3b_edge_pe(ctx, S->pe, S->delp, ptop, st));
    FV3B_CALL(fv3b_pk3_halo(ctx, pk3, S->delp, ptop, akap, st));
    // compute_geopotential (dyn_core.py:96-98) with two halo rows
    FV3B_CHECK(launch_box(Box{s - 2, e + 3, js - 2, je + 3, 0, nk}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      W3(gz, i, j) = F3(zh, i, j) * GRAV_;
    }));
    FV3B_CALL(fv3b_nh_p_grad(ctx, S->u, S->v, pkc, gz, pk3, S->delp, dt, ptop, akap, st));
    if (cfg.rf_fast)
      FV3B_CALL(fv3b_ray_fast(ctx, S->u, S->v, S->w, a->dp_ref.data(), a->pfull.data(), dt, ptop, cfg.rf_cutoff,
                              cfg.tau, 0, st));
    if (it != n_split - 1) {
      FV3B_CHECK(halo_vector(d, S->u, S->v, false, nz, st));
    } else {
      FV3B_CHECK(sync_vector_interfaces(d, S->u, S->v, nz, st));
    }
  }
  if (a->do_del2cubed) {
    FV3B_CHECK(halo_scalars(d, &heat, 1, 1, d.h, nz, st));
    FV3B_CALL(fv3b_del2cubed(ctx, heat, a->cd, dcfg.nord + 1 < 3 ? dcfg.nord + 1 : 3, st));
    const double delt_time_factor = fabs(dt * cfg.delt_max);
    FV3B_CALL(fv3b_pkz_tempadjust(ctx, S->delp, S->delz, S->cappa, heat, S->pt, S->pkz, delt_time_factor, a->nk_heat,
                                  st));
  }
  return FV3B_OK;
}

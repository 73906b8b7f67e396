// Finite-volume transport as stand-alone operators, and tracer advection.
//
// * fv3b_transport_*: FiniteVolumeTransport (fv3core/stencils/fvtp2d.py:151-362)
//   as an object, constructed with its PPM order and optional del-n damping
//   columns, called with a field and the Courant numbers and fluxes.
// * fv3b_ppm_flux: XPiecewiseParabolic / YPiecewiseParabolic
//   (xppm.py:283-347, yppm.py) over a caller-chosen box.
// * fv3b_tracer_advection: TracerAdvection (tracer_2d_1l.py:120-300), the
//   tracer transport with the acoustic loop's accumulated fluxes that
//   DynamicalCore._dyn runs after AcousticDynamics (fv_dynamics.py:544-557).
//
// All of them use the PPM and transport device code of transport.cuh, the
// same the D-grid stages use, with the ord-8 limiter for hord = 8.
#include <math.h>

#include <new>
#include <vector>

#include "halo_ops.cuh"
#include "transport.cuh"

using namespace fv3b;

namespace {

// workspace slots of these operators (none of them runs inside another
// stage); the transport's own scratch and the tracer advection's fields
constexpr int WS_TR_FX_MEAN = 33, WS_TR_FY_MEAN = 34, WS_TR_QADV_X = 35, WS_TR_QADV_Y = 36;
constexpr int WS_TR_XFX = 26, WS_TR_YFX = 27, WS_TR_FX = 28, WS_TR_FY = 29, WS_TR_DP2 = 32;
constexpr int WS_TR_DELN_FX2 = 37, WS_TR_DELN_FY2 = 38, WS_TR_DELN_D2 = 15;

bool hord_supported(int hord) { return hord == 5 || hord == 6 || hord == 7 || hord == 8; }

}  // namespace

// FiniteVolumeTransport as an object: the PPM order and, when damping is
// asked for, the per-level DelnFlux columns (calc_damp, delnflux.py:24-26,
// with da_min; the single-precision build's range scaling as in
// fv3b_d_sw_setup).
struct fv3b_transport {
  fv3b_ctx* ctx = nullptr;
  int hord = 6;
  bool damped = false;
  int nmax = 0;
  real rscale = RC(1.0);
  real* cols = nullptr;  // device [2][MAXLEV]: nord, damp
};

extern "C" int fv3b_transport_create(fv3b_ctx* ctx, int hord, const double* nord, const double* damp_c, int n,
                                     fv3b_transport** out) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && out, "fv3b_transport_create: null argument");
  FV3B_REQUIRE(hord_supported(hord), "fv3b_transport_create: hord must be 5, 6, 7 or 8");
  FV3B_REQUIRE((nord == nullptr) == (damp_c == nullptr),
               "fv3b_transport_create: give both nord and damp_c, or neither");
  const int npz = ctx->d.nz;
  fv3b_transport* tr = new (std::nothrow) fv3b_transport();
  FV3B_REQUIRE(tr != nullptr, "fv3b_transport_create: out of host memory");
  tr->ctx = ctx;
  tr->hord = hord;
  if (nord != nullptr) {
    if (n < npz || n > MAXLEV) {
      delete tr;
      FV3B_REQUIRE(false, "fv3b_transport_create: nord and damp_c need npz to 128 levels");
    }
    // DelnFlux.__init__ (delnflux.py:907-932): no damping when every
    // coefficient is small, rejected when only some below the top are
    bool all_small = true, some_small = false;
    for (int k = 0; k < n; ++k) all_small = all_small && damp_c[k] <= 1e-4;
    for (int k = 0; k < n - 1; ++k) some_small = some_small || damp_c[k] <= 1e-4;
    if (!all_small && some_small) {
      delete tr;
      set_last_error_msg("fv3b_transport_create: damp_c currently must be always greater than 10^-4 for delnflux");
      return FV3B_ERR_UNSUPPORTED;
    }
    if (!all_small) {
      double m = 0.0;
      for (int k = 0; k < n; ++k) m = nord[k] > m ? nord[k] : m;
      tr->nmax = (int)m;
      if (tr->nmax > 3) {
        delete tr;
        FV3B_REQUIRE(false, "fv3b_transport_create: nord must be less than 3");
      }
      std::vector<double> c(2 * MAXLEV, 0.0);
      for (int k = 0; k < n; ++k) c[k] = nord[k];
      for (int k = 0; k < npz; ++k) c[MAXLEV + k] = pow(damp_c[k] * ctx->m.da_min, nord[k] + 1);
      // FP32 builds: each del-n pass multiplies by a power of two near the
      // smallest area; the coefficient of a level that iterates carries
      // the inverse scale
      const bool scale_range = sizeof(real) < sizeof(double);
      const double S = scale_range ? std::ldexp(1.0, std::ilogb(ctx->m.da_min)) : 1.0;
      if (tr->nmax > 0) {
        const double f = std::pow(S, -tr->nmax);
        for (int k = 0; k < MAXLEV; ++k)
          if (c[k < 3 ? k : 3] > 0) c[MAXLEV + k] *= f;
      }
      tr->rscale = static_cast<real>(S);
      std::vector<real> cr(c.begin(), c.end());
      cudaError_t e = cudaMalloc((void**)&tr->cols, sizeof(real) * 2 * MAXLEV);
      if (e == cudaSuccess) e = cudaMemcpy(tr->cols, cr.data(), sizeof(real) * 2 * MAXLEV, cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        cudaFree(tr->cols);
        delete tr;
        set_last_error("fv3b_transport_create", e);
        return FV3B_ERR_CUDA;
      }
      tr->damped = true;
    }
  }
  *out = tr;
  return FV3B_OK;
}

extern "C" int fv3b_transport_destroy(fv3b_transport* tr) {
  if (!tr) return FV3B_OK;
  cudaError_t e = tr->cols ? cudaFree(tr->cols) : cudaSuccess;
  delete tr;
  FV3B_CHECK(e);
  return FV3B_OK;
}

namespace {

// One transport: the x corner copy of q in place on levels [0, nlev_corner),
// the three fvtp2d passes on every interface level, and the damping.
cudaError_t run_transport(const fv3b_transport* tr, real* q, const real* crx, const real* cry, const real* xfx,
                          const real* yfx, real* fx, real* fy, const real* mfx, const real* mfy, const real* mass,
                          int nlev_corner, cudaStream_t st) {
  fv3b_ctx* ctx = tr->ctx;
  const Dims d = ctx->d;
  real** W = ctx->ws;
  cudaError_t err = copy_corners_x_inplace(d, q, st, nlev_corner);
  if (err != cudaSuccess) return err;
  FvTp2dArgs a{q, crx, cry, xfx, yfx, mfx ? mfx : xfx, mfy ? mfy : yfx, fx, fy, tr->hord,
               W[WS_TR_FX_MEAN], W[WS_TR_FY_MEAN], W[WS_TR_QADV_X], W[WS_TR_QADV_Y]};
  err = fvtp2d(d, ctx->m, a, st);
  if (err != cudaSuccess || !tr->damped) return err;
  DelnCol col{tr->cols, tr->cols + MAXLEV, tr->rscale};
  return delnflux(d, ctx->m, q, fx, fy, col, mass, W[WS_TR_DELN_FX2], W[WS_TR_DELN_FY2], W[WS_TR_DELN_D2],
                  W[WS_DELN_ALT], tr->nmax, st);
}

// PPM fluxes along AXIS over a box (the body of fv3b_ppm_flux)
template <int AXIS, bool O8>
cudaError_t launch_ppm_box(const Dims d, const real* dxa, const Box b, const real* q, const real* c, real* flux,
                           int s, int e, int mord, cudaStream_t st) {
  return launch_box(b, st, [=] __device__(int t, int i, int j, int k) {
    const idx_t o = idx3(d, t, i, j, k);
    flux[o] = ppm_flux_ord<O8>(line3<AXIS>(d, q, t, i, j, k), line2<AXIS>(d, dxa, t, i, j), c[o],
                               AXIS == 0 ? i : j, s, e, mord);
  });
}

}  // namespace

extern "C" int fv3b_fvtp2d(const fv3b_transport* tr, real* q, const real* crx, const real* cry,
                           const real* x_area_flux, const real* y_area_flux, real* q_x_flux, real* q_y_flux,
                           const real* x_mass_flux, const real* y_mass_flux, const real* mass, void* stream) {
  FV3B_TILES((tr ? tr->ctx : nullptr));
  FV3B_REQUIRE(tr && q && crx && cry && x_area_flux && y_area_flux && q_x_flux && q_y_flux,
               "fv3b_fvtp2d: null argument");
  // fvtp2d.py:289-296
  FV3B_REQUIRE(!(tr->damped && mass == nullptr && (x_mass_flux != nullptr || y_mass_flux != nullptr)),
               "fv3b_fvtp2d: when damping is enabled, mass must be given if mass flux is given");
  FV3B_CHECK(run_transport(tr, q, crx, cry, x_area_flux, y_area_flux, q_x_flux, q_y_flux, x_mass_flux, y_mass_flux,
                           mass, tr->ctx->d.nk, (cudaStream_t)stream));
  return FV3B_OK;
}

// XPiecewiseParabolic.__call__ / YPiecewiseParabolic.__call__ on the box
// [i0, i0+ni) x [j0, j0+nj) x [k0, k0+nk): the mean of q advected through
// each interface of the box along the axis.
extern "C" int fv3b_ppm_flux(fv3b_ctx* ctx, int axis, int iord, const real* q, const real* c, real* flux, int i0,
                             int j0, int k0, int ni, int nj, int nk, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && q && c && flux, "fv3b_ppm_flux: null argument");
  FV3B_REQUIRE(axis == 0 || axis == 1, "fv3b_ppm_flux: axis must be 0 (x) or 1 (y)");
  FV3B_REQUIRE(hord_supported(iord), "fv3b_ppm_flux: iord must be 5, 6, 7 or 8");
  const Dims d = ctx->d;
  FV3B_REQUIRE(ni >= 0 && nj >= 0 && nk >= 0 && k0 >= 0 && k0 + nk <= d.nk, "fv3b_ppm_flux: bad vertical range");
  // the box plus the reconstruction's reach (-3..+2 along the axis) must
  // lie inside the storage
  const int lo = axis == 0 ? i0 : j0, hi = axis == 0 ? i0 + ni : j0 + nj, n_axis = axis == 0 ? d.ni : d.nj;
  const int olo = axis == 0 ? j0 : i0, ohi = axis == 0 ? j0 + nj : i0 + ni, n_other = axis == 0 ? d.nj : d.ni;
  FV3B_REQUIRE(lo - 3 >= 0 && hi + 2 <= n_axis && olo >= 0 && ohi <= n_other,
               "fv3b_ppm_flux: box and reconstruction stencil must lie inside the storage");
  if (ni == 0 || nj == 0 || nk == 0) return FV3B_OK;
  const fv3b_metrics g = ctx->m;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  const int mord = iord < 0 ? -iord : iord;
  const bool ord8 = iord == 8;
  cudaStream_t st = (cudaStream_t)stream;
  Box b{i0, i0 + ni, j0, j0 + nj, k0, k0 + nk};
  cudaError_t err;
  if (axis == 0 && ord8)
    err = launch_ppm_box<0, true>(d, g.dxa, b, q, c, flux, s, e, mord, st);
  else if (axis == 0)
    err = launch_ppm_box<0, false>(d, g.dxa, b, q, c, flux, s, e, mord, st);
  else if (ord8)
    err = launch_ppm_box<1, true>(d, g.dya, b, q, c, flux, js, je, mord, st);
  else
    err = launch_ppm_box<1, false>(d, g.dya, b, q, c, flux, js, je, mord, st);
  FV3B_CHECK(err);
  return FV3B_OK;
}

// TracerAdvection.__call__ (tracer_2d_1l.py:199-300).
extern "C" int fv3b_tracer_advection(const fv3b_transport* tr, int ntracers, real* const* tracers, real* dp1,
                                     real* mfxd, real* mfyd, real* cxd, real* cyd, double mdt, void* stream) {
  FV3B_TILES((tr ? tr->ctx : nullptr));
  (void)mdt;  // unused by the reference as well
  FV3B_REQUIRE(tr && dp1 && mfxd && mfyd && cxd && cyd && (ntracers == 0 || tracers),
               "fv3b_tracer_advection: null argument");
  FV3B_REQUIRE(ntracers >= 0, "fv3b_tracer_advection: ntracers must be >= 0");
  for (int q = 0; q < ntracers; ++q) FV3B_REQUIRE(tracers[q], "fv3b_tracer_advection: null tracer");
  fv3b_ctx* ctx = tr->ctx;
  const Dims d = ctx->d;
  const fv3b_metrics g = ctx->m;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nz = d.nz;
  cudaStream_t st = (cudaStream_t)stream;
  real** W = ctx->ws;
  real *xfx = W[WS_TR_XFX], *yfx = W[WS_TR_YFX], *fx = W[WS_TR_FX], *fy = W[WS_TR_FY];
  // flux_compute (tracer_2d_1l.py:19-60): x area flux on [is, ie+1] x
  // [js-3, je+3], y area flux on [is-3, ie+3] x [js, je+1]
  FV3B_CHECK(launch_box(Box{s - 3, e + 4, js - 3, je + 4, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    if (i >= s && i < e + 2) {
      const real cx = F3(cxd, i, j);
      W3(xfx, i, j) = cx > RC(0.0) ? cx * F2(g.dxa, i - 1, j) * F2(g.dy, i, j) * F2(g.sin_sg3, i - 1, j)
                                   : cx * F2(g.dxa, i, j) * F2(g.dy, i, j) * F2(g.sin_sg1, i, j);
    }
    if (j >= js && j < je + 2) {
      const real cy = F3(cyd, i, j);
      W3(yfx, i, j) = cy > RC(0.0) ? cy * F2(g.dya, i, j - 1) * F2(g.dx, i, j) * F2(g.sin_sg4, i, j - 1)
                                   : cy * F2(g.dya, i, j) * F2(g.dx, i, j) * F2(g.sin_sg2, i, j);
    }
  }));
  // cmax is fixed at 2 in the reference (tracer_2d_1l.py:233): 3 sub-steps,
  // and cmax_multiply_by_frac (62-81) on every storage point of npz levels
  const int n_split = (int)floor(1.0 + 2.0);
  const real frac = static_cast<real>(1.0 / n_split);
  FV3B_CHECK(launch_box(Box{0, d.ni, 0, d.nj, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    W3(cxd, i, j) = F3(cxd, i, j) * frac;
    W3(xfx, i, j) = F3(xfx, i, j) * frac;
    W3(mfxd, i, j) = F3(mfxd, i, j) * frac;
    W3(cyd, i, j) = F3(cyd, i, j) * frac;
    W3(yfx, i, j) = F3(yfx, i, j) * frac;
    W3(mfyd, i, j) = F3(mfyd, i, j) * frac;
  }));
  // the tracers' halo spec has dims (X, Y, Z): npz levels
  if (ntracers > 0) FV3B_CHECK(halo_scalars(d, tracers, ntracers, 1, d.h, nz, st));
  real *dpa = dp1, *dpb = W[WS_TR_DP2];
  for (int it = 0; it < n_split; ++it) {
    const bool last_call = it == n_split - 1;
    // dp_fluxadjustment (tracer_2d_1l.py:94-103), compute domain
    {
      const real* p1 = dpa;
      real* p2 = dpb;
      FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
        PT_SETUP(d, t, k);
        W3(p2, i, j) = F3(p1, i, j) + (F3(mfxd, i, j) - F3(mfxd, i + 1, j) + F3(mfyd, i, j) - F3(mfyd, i, j + 1)) *
                                          F2(g.rarea, i, j);
      }));
    }
    for (int q = 0; q < ntracers; ++q) {
      real* qf = tracers[q];
      // CopyCornersXY on dims (X, Y, Z): the x copy in place on npz levels
      FV3B_CHECK(run_transport(tr, qf, cxd, cyd, xfx, yfx, fx, fy, mfxd, mfyd, nullptr, nz, st));
      // q_adjust (tracer_2d_1l.py:106-128), compute domain
      const real *p1 = dpa, *p2 = dpb;
      FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
        PT_SETUP(d, t, k);
        W3(qf, i, j) = (F3(qf, i, j) * F3(p1, i, j) +
                        (F3(fx, i, j) - F3(fx, i + 1, j) + F3(fy, i, j) - F3(fy, i, j + 1)) * F2(g.rarea, i, j)) /
                       F3(p2, i, j);
      }));
    }
    if (!last_call) {
      if (ntracers > 0) FV3B_CHECK(halo_scalars(d, tracers, ntracers, 1, d.h, nz, st));
      real* tmp = dpa;
      dpa = dpb;
      dpb = tmp;
    }
  }
  return FV3B_OK;
}

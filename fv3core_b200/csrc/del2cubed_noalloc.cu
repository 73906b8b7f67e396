// fv3b_del2cubed_noalloc: the heat-source filter of HyperdiffusionDamping
// (fv3core/stencils/del2cubed.py:152-181) for callers that cannot let the
// library allocate device memory.
//
// fv3b_del2cubed takes a context, and fv3b_ctx_create allocates the whole
// stage workspace (40 full 3-D fields, tens of GB at C384) with cudaMalloc.
// Some hosts cannot allow that: a model that hands all device memory to its
// own pool (cudaMalloc from a library would fail, or fragment the pool),
// or a coupler that wants only this filter and has budgeted no memory for
// a context.  This entry point needs no context and allocates nothing.  Its
// three scratch fields live in one file-scope device array of fixed size,
// so the memory is reserved when the library's module is loaded, not when
// the call runs.
//
// Set-up: a call on a stream that is not being captured looks up the
// device address of the scratch array (cudaGetSymbolAddress, with the
// stream's device current) and keeps it per device; a call made during
// stream capture uses the kept address, so the first call on a device must
// come before any stream capture.  Looking the address up again on every
// uncaptured call keeps it valid after a cudaDeviceReset, which reloads the
// module at a new address.
//
// Sharing: there is one scratch array per device for the whole process, and
// it keeps the contents of the last call.  Nothing in it has to start at
// zero: every scratch value a call reads was written earlier in that call.
// Two calls that overlap in time on the same device (different streams, or
// different host threads without ordering) race on it and give wrong
// results.  Callers must order their calls, for example by issuing them all
// on one stream.
//
// The arithmetic is the same as fv3b_del2cubed's, launch for launch.
#include <mutex>

#include "corners.cuh"
#include "stencil.cuh"

using namespace fv3b;

namespace {

// Scratch: three fields of at most FV3B_NOALLOC_FIELD_ELEMS elements of
// fv3b_real each (6 * (npz+1) * (n+7)^2 <= 1,500,000 covers C48 L79):
// 36 MB in the FP64 build, 18 MB in the mixed-precision build.
constexpr long long FV3B_NOALLOC_FIELD_ELEMS = 1500000;
static __device__ __align__(256) real g_noalloc_scratch[3 * FV3B_NOALLOC_FIELD_ELEMS];

constexpr int MAX_DEVICES = 64;
std::mutex g_scratch_mutex;
real* g_scratch_addr[MAX_DEVICES] = {nullptr};

// Device address of the scratch array on the current device: looked up
// afresh when the stream is not capturing, the kept one otherwise.
cudaError_t scratch_address(cudaStream_t st, real** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = static_cast<real*>(p);
  } else if (g_scratch_addr[dev] == nullptr) {
    // first call on this device inside a capture: the symbol lookup may load
    // the module, which a capture does not allow
    return cudaErrorStreamCaptureUnsupported;
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int fv3b_del2cubed_noalloc(const fv3b_grid_dims* dims, const fv3b_metrics* metrics, real* qdel,
                                      double cd_in, int nmax, void* stream) {
  // the build's precision inside the kernels (the same value in FP64 builds)
  const real cd = static_cast<real>(cd_in);
  FV3B_REQUIRE(dims && metrics && qdel, "fv3b_del2cubed_noalloc: null argument");
  FV3B_REQUIRE(dims->npx >= 4 && dims->n_halo == 3 && dims->npz >= 1,
               "fv3b_del2cubed_noalloc: need npx >= 4, n_halo == 3, npz >= 1");
  FV3B_REQUIRE(dims_fit(dims), "fv3b_del2cubed_noalloc: a 3-D field of the six tiles must hold fewer than "
                               "2^31 elements");
  const Dims d = make_dims(dims);
  FV3B_REQUIRE(d.st * 6 <= FV3B_NOALLOC_FIELD_ELEMS,
               "fv3b_del2cubed_noalloc: grid too large for the static scratch "
               "(6*(npz+1)*(npx+7)^2 must be <= 1500000 elements, i.e. at most C48 L79)");
  const fv3b_metrics g = *metrics;
  real* base = nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  FV3B_CHECK(scratch_address(st, &base));
  real *q = base, *fx = base + FV3B_NOALLOC_FIELD_ELEMS, *fy = base + 2 * FV3B_NOALLOC_FIELD_ELEMS;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nz = d.nz;
  const int full = d.ni - 1;
  const int ntimes = nmax < 3 ? nmax : 3;
  for (int n = 0; n < ntimes; ++n) {
    const int nt = ntimes - (n + 1);
    // corner_fill (del2cubed.py:41-75) into q, full domain
    FV3B_CHECK(launch_box(Box{0, full, 0, full, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      const real third = RC(1.0) / RC(3.0);
      real out = F3(qdel, i, j);
      auto Q = [&](int di, int dj) { return F3(qdel, i + di, j + dj); };
      if (j == js) {
        if (i == s) out = (Q(0, 0) + Q(-1, 0) + Q(0, -1)) * third;
        else if (i == s - 1) out = (Q(1, 0) + Q(0, 0) + Q(1, -1)) * third;
        else if (i == e) out = (Q(0, 0) + Q(1, 0) + Q(0, -1)) * third;
        else if (i == e + 1) out = (Q(-1, 0) + Q(0, 0) + Q(-1, -1)) * third;
      } else if (j == js - 1) {
        if (i == s) out = (Q(0, 1) + Q(-1, 1) + Q(0, 0)) * third;
        else if (i == e) out = (Q(0, 1) + Q(1, 1) + Q(0, 0)) * third;
      } else if (j == je) {
        if (i == e) out = (Q(0, 0) + Q(1, 0) + Q(0, 1)) * third;
        else if (i == e + 1) out = (Q(-1, 0) + Q(0, 0) + Q(-1, 1)) * third;
        else if (i == s) out = (Q(0, 0) + Q(-1, 0) + Q(0, 1)) * third;
        else if (i == s - 1) out = (Q(1, 0) + Q(0, 0) + Q(1, 1)) * third;
      } else if (j == je + 1) {
        if (i == e) out = (Q(0, -1) + Q(1, -1) + Q(0, 0)) * third;
        else if (i == s) out = (Q(0, -1) + Q(-1, -1) + Q(0, 0)) * third;
      }
      W3(q, i, j) = out;
    }));
    // compute_zonal_flux / compute_meridional_flux with the corner copies of
    // q applied on read
    FV3B_CHECK(launch_box(Box{s - nt, e + 2 + nt, js - nt, je + 2 + nt, 0, nz}, st,
                          [=] __device__(int t, int i, int j, int k) {
                            PT_SETUP(d, t, k);
                            auto qx = [&](int ii, int jj) {
                              int si, sj;
                              if (nt > 0 && copy_corner_x(d, ii, jj, si, sj)) return F3(q, si, sj);
                              return F3(q, ii, jj);
                            };
                            auto qy = [&](int ii, int jj) {
                              int si, sj;
                              if (nt > 0 && copy_corner_y(d, ii, jj, si, sj)) return F3(q, si, sj);
                              return F3(q, ii, jj);
                            };
                            if (j < je + 1 + nt) W3(fx, i, j) = F2(g.del6_v, i, j) * (qx(i - 1, j) - qx(i, j));
                            if (i < e + 1 + nt) W3(fy, i, j) = F2(g.del6_u, i, j) * (qy(i, j - 1) - qy(i, j));
                          }));
    // copy back and update_q
    FV3B_CHECK(launch_box(Box{0, full, 0, full, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      int si, sj;
      real qv = (nt > 0 && copy_corner_y(d, i, j, si, sj)) ? F3(q, si, sj) : F3(q, i, j);
      if (i >= s - nt && i < e + 1 + nt && j >= js - nt && j < je + 1 + nt)
        qv = qv + cd * F2(g.rarea, i, j) * (F3(fx, i, j) - F3(fx, i + 1, j) + F3(fy, i, j) - F3(fy, i, j + 1));
      W3(qdel, i, j) = qv;
    }));
  }
  return FV3B_OK;
}

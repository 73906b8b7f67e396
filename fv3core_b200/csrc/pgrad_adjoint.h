// Hand-written adjoint (reverse mode) of p_grad_c_stencil
// (dyn_core.py:101-145, nonhydrostatic form), written for both the device
// and the host (the tests build it with g++ and compare with torch autograd
// of a PyTorch-ops restatement).
//
// The forward adds to uc and vc, at every point of [is, ie+1] x [js, je+1]
// and layer 0..npz-1, the increment
//   c * A,  c = dt2 * rdc / (delpc(q) + delpc(p)),
//   A = (gz(q, k+1) - gz(p, k)) * (pkc(p, k+1) - pkc(q, k))
//     + (gz(q, k) - gz(p, k+1)) * (pkc(q, k+1) - pkc(p, k)),
// with p the point, q its west (uc, rdc = rdxc) or south (vc, rdc = rdyc)
// neighbour.  uc and vc pass their cotangents through unchanged; the
// adjoint below gathers, for one input point, the cotangents of delpc, pkc
// and gz from the (at most eight) increments that read it, so every
// thread writes only its own point.
#pragma once

#include "dims.h"

namespace fv3b {
namespace adj {

// The terms of one increment at output offset o, neighbour o - off.
template <class R>
struct PgcTerms {
  R c, a, b, cc, e, A, D;
};

template <class R>
__host__ __device__ inline PgcTerms<R> pgc_terms(const Dims& d, const R* delpc, const R* pkc, const R* gz, R rdc,
                                                 R dt2, idx_t o, idx_t off) {
  PgcTerms<R> t;
  const idx_t q = o - off, sk = d.sk;
  t.D = delpc[q] + delpc[o];
  t.c = dt2 * rdc / t.D;
  t.a = gz[q + sk] - gz[o];
  t.b = pkc[o + sk] - pkc[q];
  t.cc = gz[q] - gz[o + sk];
  t.e = pkc[q + sk] - pkc[o];
  t.A = t.a * t.b + t.cc * t.e;
  return t;
}

// Cotangents of delpc, pkc and gz at (t, i, j, k) (k = 0..npz) from the
// cotangents gu, gv of the new uc, vc.
template <class R>
__host__ __device__ inline void pgc_point_adjoint(const Dims& d, int t, int i, int j, int k, R dt2, const R* rdxc,
                                                  const R* rdyc, const R* delpc, const R* pkc, const R* gz,
                                                  const R* gu, const R* gv, R& g_delpc, R& g_pkc, R& g_gz) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nz = d.nz;
  R a_delp = R(0), a_pk = R(0), a_gz = R(0);
  for (int face = 0; face < 2; ++face) {
    const int di = face == 0 ? 1 : 0, dj = face == 0 ? 0 : 1;
    const idx_t off = face == 0 ? 1 : d.sj;
    const R* g = face == 0 ? gu : gv;
    const R* rd = face == 0 ? rdxc : rdyc;
    // increment at (i + ei, j + ej, k + ek), ei/ej in {0, the face offset}
    auto term = [&](int ei, int ej, int ek, PgcTerms<R>& tm, R& cot) {
      const int ip = i + ei, jp = j + ej, kp = k + ek;
      if (ip < s || ip > e + 1 || jp < js || jp > je + 1 || kp < 0 || kp >= nz) return false;
      const idx_t op = idx3(d, t, ip, jp, kp);
      tm = pgc_terms<R>(d, delpc, pkc, gz, rd[idx2(d, t, ip, jp)], dt2, op, off);
      cot = g[op] * tm.c;
      return true;
    };
    PgcTerms<R> tm;
    R w;
    // the point itself as p, layer k: gz(p, k) -b, pkc(p, k) -cc, delpc(p)
    if (term(0, 0, 0, tm, w)) {
      a_gz -= w * tm.b;
      a_pk -= w * tm.cc;
      a_delp -= w * tm.A / tm.D;
    }
    // as p, layer k - 1: gz(p, k+1) -e, pkc(p, k+1) +a
    if (term(0, 0, -1, tm, w)) {
      a_gz -= w * tm.e;
      a_pk += w * tm.a;
    }
    // as q of the next point, layer k: gz(q, k) +e, pkc(q, k) -a, delpc(q)
    if (term(di, dj, 0, tm, w)) {
      a_gz += w * tm.e;
      a_pk -= w * tm.a;
      a_delp -= w * tm.A / tm.D;
    }
    // as q of the next point, layer k - 1: gz(q, k+1) +b, pkc(q, k+1) +cc
    if (term(di, dj, -1, tm, w)) {
      a_gz += w * tm.b;
      a_pk += w * tm.cc;
    }
  }
  g_delpc = k < nz ? a_delp : R(0);
  g_pkc = a_pk;
  g_gz = a_gz;
}

}  // namespace adj
}  // namespace fv3b

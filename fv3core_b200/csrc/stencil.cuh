// Point-access macros for box lambdas.  Inside a lambda called for point
// (t, i, j, k), PT_SETUP binds the tile and level; F3/W3 read/write a 3-D
// field at horizontal index (i, j) of that level, F3K at level k+dk, F2 reads
// a 2-D field of that tile.
#pragma once
#include "common.cuh"

#define PT_SETUP(d, t, k)                                  \
  const ::fv3b::idx_t _b3 = (t) * (d).st + (k) * (d).sk;   \
  const ::fv3b::idx_t _b2 = (t) * (d).st2;                 \
  const ::fv3b::idx_t _sj = (d).sj;                        \
  (void)_b3;                                               \
  (void)_b2;                                               \
  (void)_sj

#define F3(p, i, j) ((p)[_b3 + (j) * _sj + (i)])
#define W3(p, i, j) ((p)[_b3 + (j) * _sj + (i)])
#define F3K(p, i, j, dk) ((p)[_b3 + (dk) * d.sk + (j) * _sj + (i)])
#define F2(p, i, j) ((p)[_b2 + (j) * _sj + (i)])

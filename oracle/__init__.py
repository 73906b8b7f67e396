"""CPU oracle for the acoustic substep — TEST INFRASTRUCTURE ONLY.

A plain numpy FP64 restatement of the reference's (fv3core) stencils on the
acoustic-substep path.  Each function cites the reference file:line it
restates.  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg may import this package, and only as the checker or the
timed CPU baseline; the product path (``fv3core_b200``) never does.

Conventions: every function works on one cube tile; arrays are the
reference's full storages ``[n+2h+1, n+2h+1, nz+1]`` (2-D metric fields
``[n+2h+1, n+2h+1]``), indexed i, j, k.  Temporaries are evaluated over the
whole padded tile (NaN where an offset read leaves the array) and only the
reference's write domain of each output is stored, so halo contents of the
outputs match the reference exactly where it defines them.

Parity is pinned by golden fixtures produced by running the reference's own
stencil classes (``tests/golden/make_golden.py``).
"""

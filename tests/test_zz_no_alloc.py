"""fv3b_del2cubed_noalloc (no reference counterpart): the context-free,
allocation-free variant of the del2cubed filter.  It must give exactly what
fv3b_del2cubed gives, call after call, and reject grids beyond its static
scratch.  Collected last on purpose: its scratch is one fixed array shared
by the whole process."""
import ctypes

import numpy as np
import pytest

import cases
from metrics import parity_err

H = 3


def _call(name, *args):
    from fv3core_b200 import _lib

    _lib.call(name, *args)


def test_rejects_grids_beyond_the_static_scratch():
    """C64 L79 needs 6*80*71^2 = 2,419,680 elements per scratch field, over
    the 1,500,000 reserved; the call must fail before touching the device."""
    from fv3core_b200 import _lib
    from fv3core_b200.grid_data import Metrics

    dims = _lib.GridDims(64, 3, 79, 0)
    m = Metrics()
    rc = _lib.lib().fv3b_del2cubed_noalloc(ctypes.byref(dims), ctypes.addressof(m), 8, 0.1, 3, None)
    assert rc == 1  # FV3B_ERR_ARGUMENT
    assert b"static scratch" in _lib.lib().fv3b_last_error()


def test_rejects_grids_beyond_32_bit_offsets_with_their_own_message():
    from fv3core_b200 import _lib
    from fv3core_b200.grid_data import Metrics

    dims = _lib.GridDims(2000, 3, 150, 0)
    m = Metrics()
    rc = _lib.lib().fv3b_del2cubed_noalloc(ctypes.byref(dims), ctypes.addressof(m), 8, 0.1, 3, None)
    assert rc == 1  # FV3B_ERR_ARGUMENT
    assert b"2^31" in _lib.lib().fv3b_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("n,nz,precision", [(12, 8, "f64"), (48, 79, "f64"), (12, 8, "f32"), (48, 79, "f32")])
def test_matches_context_entry_point_on_consecutive_calls(n, nz, precision):
    """Both builds: the FP64 library to the last bit; the mixed-precision
    library (its own fixed scratch of FP32 elements) within a few FP32 ulps
    (1e-6 relative), since that build lets the compiler contract a*b+c in
    each kernel on its own."""
    import torch

    from fv3core_b200 import _lib
    from fv3core_b200.grid_data import GridData
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils.del2cubed import HyperdiffusionDamping
    from fv3core_b200.storage import stream_ptr, to_device, to_host

    gd = GridData(cases.grid_for(n), nz, precision=precision)
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    dtype = gd.grid_indexing.dtype
    rng = np.random.default_rng(n + nz)
    m = n + 2 * H + 1
    g = cases.grid_for(n)
    cd = 0.2 * g.da_min
    damp = HyperdiffusionDamping(sf, gd, gd.rarea, 3)
    dims = gd.grid_indexing.dims()
    try:
        for call in range(2):
            heat = 1e3 * rng.standard_normal((6, m, m, nz + 1))
            a, b = to_device(heat, dtype=dtype), to_device(heat, dtype=dtype)
            damp(a, cd)
            _lib.call("fv3b_del2cubed_noalloc", dims, ctypes.addressof(gd._metrics), b.data_ptr(), cd, 3,
                      stream_ptr(), precision=precision)
            torch.cuda.synchronize()
            if precision == "f64":
                assert np.array_equal(to_host(a), to_host(b)), call
            else:
                assert parity_err(to_host(b), to_host(a)) <= 1e-6, call
    finally:
        gd.close()
